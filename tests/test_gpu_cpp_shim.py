"""The C++ classes of include/wahgpu.hpp (bitvector, relic, bin,
countQuery with WHERE clauses), compiled with g++ and run on the GPU, give
the reference's words and the scans' row sets."""
import os
import struct
import subprocess
import tempfile

import numpy as np
import pytest

from conftest import load_golden, unpack
from test_gpu_build import canonical_words
import oracle
from oracle import wahgen as G

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _build(td):
    exe = os.path.join(td, "shim_test")
    cuda = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    lib = os.path.join(ROOT, "libfastlib_b200")
    subprocess.run(["g++", "-std=c++17", "-O1", "-I" + os.path.join(ROOT, "include"), "-I" + cuda + "/include",
                    os.path.join(ROOT, "tests", "cpp", "shim_test.cpp"), "-o", exe,
                    "-L" + lib, "-lwahgpu", "-Wl,-rpath," + lib, "-L" + cuda + "/lib64", "-lcudart"],
                   check=True)
    return exe


def _u32v(a):
    a = np.asarray(a, dtype=np.uint32)
    return struct.pack("<I", len(a)) + a.tobytes()


class _R:
    def __init__(self, data):
        self.d, self.p = data, 0

    def u64(self):
        v = struct.unpack_from("<Q", self.d, self.p)[0]
        self.p += 8
        return v

    def vec(self):
        n = self.u64()
        v = np.frombuffer(self.d, np.uint32, n, self.p).copy()
        self.p += 4 * n
        return v


def test_cpp_shim(gpu_ctx):
    g = load_golden("binop_random.npz")
    cases = []
    for i in range(len(g["op"])):
        if g["status"][i] != 0 or len(cases) >= 120:
            continue
        a, b = unpack(g, "a", i), unpack(g, "b", i)
        if oracle.is_degenerate(a) or oracle.is_degenerate(b):
            continue
        cases.append((int(g["op"][i]), int(g["inplace"][i]), a, b, unpack(g, "res", i), int(g["cnt"][i])))
    rng = np.random.default_rng(3)
    builds = []
    for nbits in (1, 40, 62, 1000, 5000):
        rows = np.unique(rng.integers(0, nbits, max(1, nbits // 7)))
        if nbits >= 1000:
            rows = np.unique(np.concatenate([rows, np.arange(100, 200)]))  # all-1 groups
        builds.append((nbits, rows.astype(np.uint32)))
    n = 100_003
    ca = rng.integers(0, 100, n).astype(np.uint32)
    cb = rng.normal(0, 1, n).astype(np.float32)
    clauses = ["a >= 10 and a < 20", "a between 5 and 7 and b < 0.5", "0.25 <= b < 1.5", "b > -0.3 and a = 42",
               "A <= 3", "a < 50 and b >= 0 and a > 40", "c < 3", "a < 5 or b < -1", "not a < 50",
               "a != 42 and b < 0", "(a < 10 or a >= 90) and not (b between -0.5 and 0.5)", "!(a >= 3) || b > 2",
               "a < 5 or", "(a < 3", "a < 20 and (b < -1 or b > 1) and a >= 10", "a in (3, 17, 42) or b > 2.5",
               "a in (3, 17"]
    data = struct.pack("<I", len(cases))
    for op, ip, a, b, _, _ in cases:
        data += struct.pack("<II", op, ip) + _u32v(a) + _u32v(b)
    data += struct.pack("<I", len(builds))
    for nbits, rows in builds:
        data += struct.pack("<I", nbits) + _u32v(rows)
    data += struct.pack("<I", n) + _u32v(ca) + _u32v(cb.view(np.uint32))
    data += struct.pack("<I", len(clauses))
    for c in clauses:
        data += _u32v([ord(ch) for ch in c])
    # section 5: array-like constructor, setBit inside, shrinking adjustSize
    arr = oracle.build_runs(G.geometric_runs(31, 20000, 0.2))
    arr_bits = np.zeros(20000, bool)
    arr_bits[oracle.rids(arr)] = True
    set_at = int(np.flatnonzero(~arr_bits)[100])
    clear_at = int(np.flatnonzero(arr_bits)[50])
    keep = 12345
    data += _u32v(arr) + struct.pack("<III", set_at, clear_at, keep)
    with tempfile.TemporaryDirectory() as td:
        exe = _build(td)
        fi, fo = os.path.join(td, "in.bin"), os.path.join(td, "out.bin")
        open(fi, "wb").write(data)
        gold = os.path.join(ROOT, "tests", "golden")
        subprocess.run([exe, fi, fo, os.path.join(gold, "relic_3001.idx"), os.path.join(gold, "bin_5000.idx")],
                       check=True)
        R = _R(open(fo, "rb").read())
    for k, (op, ip, a, b, res, cnt) in enumerate(cases):
        assert np.array_equal(R.vec(), res), k
        assert R.u64() == cnt, k
    for nbits, rows in builds:
        assert np.array_equal(R.vec(), canonical_words(rows, nbits)), nbits
        assert np.array_equal(R.vec(), rows), nbits
        assert np.array_equal(R.vec(), canonical_words(rows, nbits + 45)), nbits
        assert R.u64() == len(rows), nbits
    fa, fb = ca.astype(np.float64), cb.astype(np.float64)
    want = [(fa >= 10) & (fa < 20), (fa >= 5) & (fa <= 7) & (fb < 0.5), (fb >= 0.25) & (fb < 1.5),
            (fb > -0.3) & (fa == 42), fa <= 3, (fa < 50) & (fb >= 0) & (fa > 40), None, (fa < 5) | (fb < -1),
            ~(fa < 50), (fa != 42) & (fb < 0), ((fa < 10) | (fa >= 90)) & ~((fb >= -0.5) & (fb <= 0.5)),
            ~(fa >= 3) | (fb > 2), None, None, (fa < 20) & ((fb < -1) | (fb > 1)) & (fa >= 10),
            np.isin(fa, [3, 17, 42]) | (fb > 2.5), None]
    for c, m in zip(clauses, want):
        rc = struct.unpack("<q", struct.pack("<Q", R.u64()))[0]
        if m is None:
            assert rc < 0, c
            continue
        assert rc == 0, c
        assert R.u64() == m.sum(), c
        assert np.array_equal(R.vec(), np.flatnonzero(m)), c
    m = (fa >= 10) & (fa < 20)
    assert R.u64() == m.sum() and R.u64() == m.sum()
    assert np.array_equal(R.vec(), np.flatnonzero(m))
    # bin estimate: lower holds only hits, upper (or lower when upper is
    # empty) holds every hit, and the count bound covers it
    hits = set(np.flatnonzero((fb >= -0.5) & (fb < 0.25)).tolist())
    lower = R.vec()
    usize = R.u64()
    upper = R.vec()
    bound = R.u64()
    assert set(lower.tolist()) <= hits
    sup = set(upper.tolist()) if usize else set(lower.tolist())
    assert hits <= sup and bound == len(sup)
    # relic read from the reference-written file; a bin file refused as relic
    rv = load_golden("idxfile_inputs.npz")["relic_vals"].astype(np.float64)
    m = (rv >= 10) & (rv < 30)
    assert R.u64() == m.sum()
    assert np.array_equal(R.vec(), np.flatnonzero(m))
    assert R.u64() == 1
    # array-like constructor, setBit inside the vector, shrinking adjustSize
    bits = arr_bits.copy()
    bits[set_at] = True
    bits[clear_at] = False
    assert np.array_equal(R.vec(), np.flatnonzero(bits))
    assert R.u64() == keep
    assert np.array_equal(R.vec(), np.flatnonzero(bits[:keep]))
