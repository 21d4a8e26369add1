"""Host-only parts of the C++ classes (include/wahgpu.hpp), compiled with
g++ and run without a device: the indexSet walk (src/bitvector.h:421-522,
src/bitvector.cpp:4524-4590) yields the oracle's row ids for the golden
operands and generated word forms, and the truncation of a shrinking
adjustSize (erase, src/bitvector.cpp:1012-1036) keeps exactly the first nt
bits in a valid serialized form."""
import os
import struct
import subprocess
import tempfile

import numpy as np
import pytest

import oracle
from oracle import wahgen as G
from conftest import load_golden, unpack

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "libfastlib_b200")


@pytest.fixture(scope="module")
def exe():
    if not os.path.exists(os.path.join(LIB, "libwahgpu.so")):
        pytest.skip("libwahgpu.so not built")
    td = tempfile.mkdtemp()
    out = os.path.join(td, "host_shim_test")
    cuda = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    subprocess.run(["g++", "-std=c++17", "-O1", "-I" + os.path.join(ROOT, "include"), "-I" + cuda + "/include",
                    os.path.join(ROOT, "tests", "cpp", "host_shim_test.cpp"), "-o", out,
                    "-L" + LIB, "-lwahgpu", "-Wl,-rpath," + LIB, "-L" + cuda + "/lib64", "-lcudart"], check=True)
    return out


def _cases():
    g = load_golden("binop_random.npz")
    cases = [unpack(g, "a", i) for i in range(0, len(g["op"]), 7)]
    rng = np.random.default_rng(9)
    for style in ("mixed", "short", "dense", "sparse", "canon"):
        for _ in range(6):
            ng = int(rng.integers(0, 300))
            cases.append(np.asarray(G.serialize(G.random_words(rng, ng, style), int(rng.integers(0, 31)),
                                                int(rng.integers(0, 1 << 31))), np.uint32))
    cases.append(np.asarray([0], np.uint32))               # empty
    cases.append(np.asarray([0x15, 5], np.uint32))         # active word only
    return cases


def _bits(ser):
    """Bit array of a serialized bitvector (row order)."""
    ser = np.asarray(ser, np.uint32)
    n = oracle._groups(ser) * 31 + (int(ser[-1]) if 0 < ser[-1] < 31 else 0)
    b = np.zeros(n, bool)
    b[oracle.rids(ser)] = True
    return b


def test_index_set_and_truncate(exe):
    cases = _cases()
    rng = np.random.default_rng(10)
    keeps = []
    for ser in cases:
        n = len(_bits(ser))
        keeps.append(int(rng.integers(0, n + 1)) if n else 0)
    req = struct.pack("<I", len(cases)) + b"".join(
        struct.pack("<II", k, len(s)) + np.asarray(s, np.uint32).tobytes() for s, k in zip(cases, keeps))
    with tempfile.TemporaryDirectory() as td:
        fi, fo = os.path.join(td, "in"), os.path.join(td, "out")
        open(fi, "wb").write(req)
        subprocess.run([exe, fi, fo], check=True)
        d = open(fo, "rb").read()
    p = 0
    for ser, keep in zip(cases, keeps):
        n = struct.unpack_from("<I", d, p)[0]
        pos = np.frombuffer(d, np.uint32, n, p + 4)
        p += 4 + 4 * n
        assert np.array_equal(pos, oracle.rids(ser))
        n = struct.unpack_from("<I", d, p)[0]
        t = np.frombuffer(d, np.uint32, n, p + 4)
        p += 4 + 4 * n
        tb = _bits(t)
        assert len(tb) == keep
        assert np.array_equal(tb, _bits(ser)[:keep])
